"""Host mirror of the legacy dry preheat over the CUDA kernels.

`Preheat` keeps the shape of mantle::couple::AdvanceLegacyPreheat
(src/couple/preheat.h:26, preheat.cpp:235-287): H advected by the frozen
Stokes velocity and diffused, C fixed, forward Euler with a step bounded by
cfl / the constant per-cell rate of Build (preheat.cpp:65-159). `run()` is
AdvanceLegacyPreheat (history rows as PreheatStep, a PreheatReport, and the
diagnostic T and phi); `begin`/`advance`/`rhs`/`diagnostics` expose its parts.
`write_history` writes preheat_history.csv as WritePreheatHistory
(preheat.cpp:289-312). Arrays may be numpy (host) or CUDA tensors.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np
import torch

from . import _capi
from .synthetic import Material, Workload, material_s

STEP_FIELDS = [n for n, _ in _capi.PreheatStep._fields_]
REPORT_FIELDS = [n for n, _ in _capi.PreheatReport._fields_]
HISTORY_COLUMNS = "step,time,time_years,dt,dt_s,courant,H_integral,h_mean_J_kg,h_min_J_kg,h_max_J_kg,outward_H_flux,balance_error"


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        return a.data_ptr()
    return a.ctypes.data


def _host(a):
    if isinstance(a, torch.Tensor):
        return a
    return np.ascontiguousarray(a, dtype=np.float64)


def _row(r) -> dict:
    return {n: getattr(r, n) for n in STEP_FIELDS}


@dataclasses.dataclass
class PreheatConfig:
    """The Configuration subset the preheat reads (input time controls,
    transport boundary rules, stabilizer, thermal diffusivity, phase model)."""
    material: Material = dataclasses.field(default_factory=material_s)
    pressure_model: int = 0          # 0 constant (pressure Pa), 1 lithostatic (pressure = surface_y)
    pressure: float = 0.0
    end: float = 1.0
    max_steps: int = 100000
    control: int = 0                 # 0 cfl, 1 fixed
    dt_initial: float = 1e-3
    dt_min: float = 1e-8
    dt_max: float = 1e-2
    cfl: float = 0.5
    diffusivity: float = 0.0
    thermal_type: tuple = (0, 0, 0, 0)       # walls bottom, top, left, right
    thermal_value: tuple = (0.0, 0.0, 0.0, 0.0)
    H_policy: int = 0
    inflow_H: float = 1.0
    lf_global: int = 0
    lf_global_speed: float = 0.0

    def to_c(self) -> _capi.PreheatOpts:
        m = _capi.Material(*[float(x) for x in dataclasses.astuple(self.material)])
        return _capi.PreheatOpts(m, int(self.pressure_model), float(self.pressure), float(self.end),
                                 int(self.max_steps), int(self.control), float(self.dt_initial),
                                 float(self.dt_min), float(self.dt_max), float(self.cfl), float(self.diffusivity),
                                 (C.c_int * 4)(*[int(x) for x in self.thermal_type]),
                                 (C.c_double * 4)(*[float(x) for x in self.thermal_value]),
                                 int(self.H_policy), float(self.inflow_H), int(self.lf_global),
                                 float(self.lf_global_speed))


class Preheat:
    """One preheat instance resident on the GPU."""

    CFL, FIXED = 0, 1

    def __init__(self, w: Workload, config: PreheatConfig | None = None, stream=None, vertices=None):
        """vertices: (nx+1)*(ny+1) (x, y) pairs of a general quad mesh
        (mp_preheat_create_quads); None for the uniform mesh of w."""
        self._lib = _capi.lib()
        self.w = w
        self.config = config or PreheatConfig()
        mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
        opts = self.config.to_c()
        h = C.c_void_p()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        if vertices is None:
            _capi.check(self._lib.mp_preheat_create(C.byref(mesh), C.byref(opts), s, C.byref(h)))
        else:
            xy = np.ascontiguousarray(vertices, dtype=np.float64)
            _capi.check(self._lib.mp_preheat_create_quads(C.byref(mesh), xy.ctypes.data, C.byref(opts), s,
                                                           C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mp_preheat_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_velocity(self, vn):
        """Normal Stokes velocity at the edge Gauss points, [edge*5 + q]."""
        v = _host(vn)
        _capi.check(self._lib.mp_preheat_set_velocity(self._h, _ptr(v)))

    def set_state(self, H, Cc, time: float = 0.0, accepted: int = 0):
        Hh, Ch = _host(H), _host(Cc)
        _capi.check(self._lib.mp_preheat_set_state(self._h, _ptr(Hh), _ptr(Ch), float(time), int(accepted)))

    def get_state(self):
        H = np.zeros(self.w.cells)
        t, a = C.c_double(), C.c_longlong()
        _capi.check(self._lib.mp_preheat_get_state(self._h, _ptr(H), C.byref(t), C.byref(a)))
        return H, t.value, a.value

    def get_state_into(self, H):
        t, a = C.c_double(), C.c_longlong()
        _capi.check(self._lib.mp_preheat_get_state(self._h, _ptr(H), C.byref(t), C.byref(a)))
        return t.value, a.value

    def begin(self):
        """Build: (per-cell rate, step limit, first history row)."""
        rate = np.zeros(self.w.cells)
        limit = C.c_double()
        first = _capi.PreheatStep()
        _capi.check(self._lib.mp_preheat_begin(self._h, _ptr(rate), C.byref(limit), C.byref(first)))
        return rate, limit.value, _row(first)

    def rhs(self):
        """(dH/dt, outward boundary flux) of the current H."""
        r = np.zeros(self.w.cells)
        b = C.c_double()
        _capi.check(self._lib.mp_preheat_rhs(self._h, _ptr(r), C.byref(b)))
        return r, b.value

    def advance(self, nsteps: int, raise_on_error: bool = True):
        """Up to nsteps steps; returns (status, rows)."""
        rows = (_capi.PreheatStep * max(1, nsteps))()
        taken = C.c_longlong()
        code = self._lib.mp_preheat_advance(self._h, C.c_longlong(nsteps), rows, C.byref(taken))
        if code and raise_on_error:
            _capi.check(code)
        return code, [_row(r) for r in rows[:taken.value]]

    def diagnostics(self):
        T, phi = np.zeros(self.w.cells), np.zeros(self.w.cells)
        _capi.check(self._lib.mp_preheat_diagnostics(self._h, _ptr(T), _ptr(phi)))
        return T, phi

    def run(self, capacity: int = 100000, raise_on_error: bool = True):
        """AdvanceLegacyPreheat: (status, report, history rows, T, phi)."""
        hist = (_capi.PreheatStep * max(1, capacity))()
        rep = _capi.PreheatReport()
        n = C.c_longlong()
        T, phi = np.zeros(self.w.cells), np.zeros(self.w.cells)
        code = self._lib.mp_preheat_run(self._h, C.byref(rep), hist, C.c_longlong(capacity), C.byref(n),
                                        _ptr(T), _ptr(phi))
        if code and raise_on_error:
            _capi.check(code)
        rows = [_row(r) for r in hist[:min(n.value, capacity)]]
        return code, {k: getattr(rep, k) for k in REPORT_FIELDS}, rows, T, phi


def write_history(path: str, rows: list[dict], derived: dict, domain: tuple[float, float, float, float]) -> None:
    """preheat_history.csv with the reference's columns and 17 significant
    digits (WritePreheatHistory, preheat.cpp:289-312); written to a temporary
    name and renamed."""
    x0, x1, y0, y1 = domain
    area = (x1 - x0) * (y1 - y0)
    year = 365 * 24 * 3600
    g = lambda v: format(float(v), ".17g")
    lines = [HISTORY_COLUMNS]
    for r in rows:
        vals = [r["time"], r["time"] * derived["t0"] / year, r["dt"], r["dt"] * derived["t0"], r["courant"],
                r["integral"], r["integral"] / area * derived["h0"], r["minimum"] * derived["h0"],
                r["maximum"] * derived["h0"], r["boundaryFlux"], r["balanceError"]]
        lines.append(f"{int(r['step'])}," + ",".join(g(v) for v in vals))
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(lines) + "\n")
    os.replace(tmp, path)

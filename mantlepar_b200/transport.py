"""Host mirror of the coupled H/C transport step over the CUDA kernels.

`Transport` keeps the shape of mantle::couple::AdvancePhaseCoupled
(src/couple/evolve.h:17) and its stage RHS (src/couple/evolve.cpp:279):
create from a mesh + configuration subset, load the flow supplier's face
velocities and a cell-average state, then `rhs()` for one stage or
`step(n)` for n accepted steps of the CFL-controlled SSP Runge-Kutta loop.
Arrays may be numpy (host) or CUDA tensors; the kernels always run on the GPU.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np
import torch

from . import _capi
from .synthetic import Material, Workload, material_s

REPORT_FIELDS = [n for n, _ in _capi.StepReport._fields_]


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        return a.data_ptr()
    return a.ctypes.data


def _host(a) -> np.ndarray:
    if isinstance(a, torch.Tensor):
        return a
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclasses.dataclass
class TransportConfig:
    material: Material = dataclasses.field(default_factory=material_s)
    pressure: float = 0.0
    cfl: float = 0.4
    dt_initial: float = 1e30
    dt_max: float = 1e30
    dt_min: float = 1e-14
    theta: float = 0.0
    inflow_H: float = 1.0
    inflow_C: float = 0.3
    H_policy: int = 0
    C_policy: int = 0
    integrator: int = 3
    lf_global: int = 0
    lf_global_speed: float = 0.0
    diffusivity: float = 0.0
    precision: int = 0

    def to_c(self) -> _capi.TransportOpts:
        m = _capi.Material(*[float(x) for x in dataclasses.astuple(self.material)])
        return _capi.TransportOpts(m, self.pressure, self.cfl, self.dt_initial, self.dt_max, self.dt_min,
                                   self.theta, self.inflow_H, self.inflow_C, self.H_policy, self.C_policy,
                                   self.integrator, self.lf_global, self.lf_global_speed, self.diffusivity,
                                   self.precision)


class Transport:
    """One transport instance resident on the GPU."""

    def __init__(self, w: Workload, config: TransportConfig | None = None, stream=None, vertices=None):
        """vertices: (nx+1)*(ny+1) (x, y) pairs of a general quad mesh
        (mp_transport_create_quads); None for the uniform mesh of w."""
        self._lib = _capi.lib()
        self.w = w
        self.config = config or TransportConfig(cfl=w.cfl, integrator=w.integrator)
        mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
        opts = self.config.to_c()
        h = C.c_void_p()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        if vertices is None:
            _capi.check(self._lib.mp_transport_create(C.byref(mesh), C.byref(opts), s, C.byref(h)))
        else:
            xy = np.ascontiguousarray(vertices, dtype=np.float64)
            _capi.check(self._lib.mp_transport_create_quads(C.byref(mesh), xy.ctypes.data, C.byref(opts), s,
                                                             C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mp_transport_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_face_velocity(self, vs_n, ud_n):
        vs, ud = _host(vs_n), _host(ud_n)
        _capi.check(self._lib.mp_transport_set_face_velocity(self._h, _ptr(vs), _ptr(ud)))

    def set_state(self, H, Cc, time: float = 0.0):
        Hh, Ch = _host(H), _host(Cc)
        _capi.check(self._lib.mp_transport_set_state(self._h, _ptr(Hh), _ptr(Ch), float(time)))

    def get_state(self):
        n = self.w.cells
        H, Cc, T, phi = (np.zeros(n) for _ in range(4))
        _capi.check(self._lib.mp_transport_get_state(self._h, _ptr(H), _ptr(Cc), _ptr(T), _ptr(phi)))
        return H, Cc, T, phi

    def get_state_into(self, H=None, Cc=None, T=None, phi=None):
        _capi.check(self._lib.mp_transport_get_state(self._h, _ptr(H), _ptr(Cc), _ptr(T), _ptr(phi)))

    def rhs(self):
        n = self.w.cells
        rh, rc, T, phi, rate = (np.zeros(n) for _ in range(5))
        tot = _capi.StageTotals()
        _capi.check(self._lib.mp_transport_rhs(self._h, _ptr(rh), _ptr(rc), _ptr(T), _ptr(phi), _ptr(rate), C.byref(tot)))
        return dict(rhsH=rh, rhsC=rc, T=T, phi=phi, rate=rate,
                    **{k: getattr(tot, k) for k, _ in _capi.StageTotals._fields_})

    def limiter(self):
        n = self.w.cells
        a, b = np.zeros(n), np.zeros(n)
        _capi.check(self._lib.mp_transport_limiter(self._h, _ptr(a), _ptr(b)))
        return a, b

    CFL, FIXED = 0, 1
    ZERO_FLUX, TEMPERATURE, FLUX = 0, 1, 2

    CONSTANT, LITHOSTATIC = 0, 1

    def set_pressure_model(self, model: int, value: float):
        """CONSTANT (value: pressure in Pa) or LITHOSTATIC (value: surface_y)."""
        _capi.check(self._lib.mp_transport_set_pressure_model(self._h, int(model), float(value)))

    def set_cell_velocity(self, vs_y, ud_y):
        """Vertical solid / Darcy velocity at the cell quadrature points [cell*25 + b*5 + a]."""
        a, b = _host(vs_y), _host(ud_y)
        _capi.check(self._lib.mp_transport_set_cell_velocity(self._h, _ptr(a), _ptr(b)))

    def set_thermal_bc(self, types=(0, 0, 0, 0), values=(0.0, 0.0, 0.0, 0.0)):
        """Thermal conditions per wall (bottom, top, left, right): ZERO_FLUX,
        TEMPERATURE (dimensionless T) or FLUX (outward diffusive flux per length)."""
        ti = (C.c_int * 4)(*[int(x) for x in types])
        tv = (C.c_double * 4)(*[float(x) for x in values])
        _capi.check(self._lib.mp_transport_set_thermal_bc(self._h, ti, tv))

    def set_time_control(self, control: int, t_end: float = float("inf")):
        """time.control ("cfl" = CFL, "fixed" = FIXED) and time.end of the coupled loop."""
        _capi.check(self._lib.mp_transport_set_time_control(self._h, int(control), float(t_end)))

    def get_time(self):
        t, n = C.c_double(0.0), C.c_int(0)
        _capi.check(self._lib.mp_transport_get_time(self._h, C.byref(t), C.byref(n)))
        return t.value, n.value

    def step(self, nsteps: int, raise_on_error: bool = True):
        reps = (_capi.StepReport * max(1, nsteps))()
        code = self._lib.mp_transport_step(self._h, int(nsteps), reps)
        out = [{k: getattr(r, k) for k in REPORT_FIELDS} for r in reps[:nsteps]]
        if raise_on_error:
            _capi.check(code)
        return code, out


    def set_device_steps(self, enable: bool = True):
        """step() as CUDA graphs with the step decisions on the device (default)
        or as the host-driven loop (one device->host read per stage)."""
        _capi.check(self._lib.mp_transport_set_device_steps(self._h, int(enable)))

    def host_syncs(self) -> int:
        """Host waits for device results made by step() and rhs() so far."""
        n = C.c_ulonglong(0)
        _capi.check(self._lib.mp_transport_run_stats(self._h, C.byref(n)))
        return n.value

    def profile(self, enable: bool = True):
        """Per-kernel CUDA-event timing on (resets the accumulators) or off."""
        _capi.check(self._lib.mp_transport_profile(self._h, int(enable)))

    def kernel_times(self):
        """(ms[6], launches[6]) accumulated since profile(True): reconstruction
        (on a general quad mesh: the whole reconstruction, cell phase and face
        work), cell phase, faces, accumulation, axpy and reductions."""
        ms = (C.c_double * 6)()
        n = (C.c_ulonglong * 6)()
        _capi.check(self._lib.mp_transport_kernel_times(self._h, ms, n))
        return list(ms), list(n)


def mesh_vertices(w: Workload, family: int, perturbation: float = 0.0, seed: int = 1) -> np.ndarray:
    """Vertices of a reference mesh family from the library (mp_mesh_vertices)."""
    xy = np.zeros(2 * (w.nx + 1) * (w.ny + 1))
    mesh = _capi.MeshDesc(w.nx, w.ny, w.x0, w.x1, w.y0, w.y1)
    _capi.check(_capi.lib().mp_mesh_vertices(C.byref(mesh), int(family), float(perturbation), int(seed),
                                             xy.ctypes.data))
    return xy

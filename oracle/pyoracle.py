"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (the restatement) and, where it was built,
``oracle/_ref/libmpref.so`` (the reference's own sources compiled with the
serial stand-ins).  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline legs import this module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
FP64_PATH = os.path.join(HERE, "liboracle_fp64.so")
REF_PATH = os.path.join(HERE, "_ref", "libmpref.so")

PHASE_FIELDS = ["phi1", "phi2", "phil", "cl", "cs", "region", "TDp", "Tep",
                "dTD_dCD", "dTD_dHD", "has_solid", "has_liquid",
                "finite_temperature_derivatives"]


class Material(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ["Tm0", "Te0", "nu", "L", "cp", "Xe", "rho", "rhor", "mus", "mul", "k0", "g", "alpha0"]]


class Derived(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ["dT", "h0", "gamma", "LD", "TDm0", "TDe0", "invk0", "l0", "u0", "p0", "t0"]]


class Bounds(C.Structure):
    _fields_ = [(n, C.c_double) for n in ["Tep", "Tmp", "H_eutectic_end", "H_liquidus"]]


class Phase(C.Structure):
    _fields_ = [("phi1", C.c_double), ("phi2", C.c_double), ("phil", C.c_double),
                ("cl", C.c_double), ("cs", C.c_double), ("region", C.c_int),
                ("TDp", C.c_double), ("Tep", C.c_double), ("dTD_dCD", C.c_double),
                ("dTD_dHD", C.c_double), ("has_solid", C.c_int), ("has_liquid", C.c_int),
                ("finite_temperature_derivatives", C.c_int)]


PHASE_DTYPE = np.dtype([("phi1", "f8"), ("phi2", "f8"), ("phil", "f8"), ("cl", "f8"), ("cs", "f8"),
                        ("region", "i4"), ("TDp", "f8"), ("Tep", "f8"), ("dTD_dCD", "f8"),
                        ("dTD_dHD", "f8"), ("has_solid", "i4"), ("has_liquid", "i4"),
                        ("finite_temperature_derivatives", "i4")], align=True)
assert PHASE_DTYPE.itemsize == C.sizeof(Phase)


class TransportOpts(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("x0", C.c_double), ("x1", C.c_double),
                ("y0", C.c_double), ("y1", C.c_double), ("pressure", C.c_double), ("cfl", C.c_double),
                ("dt_initial", C.c_double), ("dt_max", C.c_double), ("dt_min", C.c_double),
                ("theta", C.c_double), ("inflow_H", C.c_double), ("inflow_C", C.c_double),
                ("H_policy", C.c_int), ("C_policy", C.c_int), ("integrator", C.c_int),
                ("lf_global", C.c_int), ("lf_global_speed", C.c_double),
                ("uniform_tables", C.c_int), ("threads", C.c_int), ("mesh_family", C.c_int),
                ("perturbation", C.c_double), ("seed", C.c_ulonglong)]


class StepReport(C.Structure):
    _fields_ = [("status", C.c_int), ("retries", C.c_int), ("dt", C.c_double), ("time", C.c_double),
                ("courant", C.c_double), ("boundaryH", C.c_double), ("boundaryC", C.c_double),
                ("sourceH", C.c_double), ("maxRate", C.c_double), ("divergence", C.c_double),
                ("balanceH", C.c_double), ("balanceC", C.c_double), ("H_integral", C.c_double),
                ("C_integral", C.c_double)]


class PreheatStep(C.Structure):
    _fields_ = [("step", C.c_longlong), ("time", C.c_double), ("dt", C.c_double), ("courant", C.c_double),
                ("integral", C.c_double), ("minimum", C.c_double), ("maximum", C.c_double),
                ("boundaryFlux", C.c_double), ("balanceError", C.c_double)]


def _row(r) -> dict:
    return {n: getattr(r, n) for n, _ in PreheatStep._fields_}


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


class _Lib:
    def __init__(self, path: str, prefix: str):
        self.lib = C.CDLL(path)
        self.prefix = prefix
        L = self.lib
        for name in ["phase_derive", "phase_boundaries", "phase_evaluate", "phase_classify",
                     "phase_evaluate_batch"]:
            getattr(L, f"{prefix}_{name}").restype = C.c_int
        t = lambda n: getattr(L, f"{prefix}_transport_{n}")
        t("create").restype = C.c_void_p
        t("create").argtypes = [C.POINTER(Material), C.POINTER(TransportOpts)]
        t("destroy").argtypes = [C.c_void_p]
        for n in ["set_face_velocity", "set_state", "get_state", "rhs", "limiter", "step", "set_time_control",
                  "set_diffusion", "set_pressure_model", "set_cell_velocity"]:
            t(n).restype = C.c_int
        t("set_pressure_model").argtypes = [C.c_void_p, C.c_int, C.c_double]
        t("set_cell_velocity").argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        t("set_diffusion").argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        t("set_time_control").argtypes = [C.c_void_p, C.c_int, C.c_double]
        t("set_face_velocity").argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        t("set_state").argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double]
        t("get_state").argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 4
        t("rhs").argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 5 + [C.POINTER(StepReport)]
        t("limiter").argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        t("step").argtypes = [C.c_void_p, C.c_int, C.POINTER(StepReport)]
        t("vertices").restype = C.c_int
        t("vertices").argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        p = lambda n: getattr(L, f"{prefix}_preheat_{n}")
        for n in ["begin", "rhs", "advance", "diagnostics"]:
            p(n).restype = C.c_int
        p("begin").argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(PreheatStep)]
        p("rhs").argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        p("advance").argtypes = [C.c_void_p, C.c_longlong, C.c_longlong, C.POINTER(PreheatStep),
                                 C.POINTER(C.c_longlong)]
        p("diagnostics").argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]

    def f(self, name):
        return getattr(self.lib, f"{self.prefix}_{name}")


_LIBS: dict[str, _Lib] = {}


def restated() -> "_Lib":
    if "orc" not in _LIBS:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        _LIBS["orc"] = _Lib(LIB_PATH, "orc")
    return _LIBS["orc"]


def restated_fp64() -> "_Lib":
    """The restatement with its per-cell and per-face steps in double instead
    of the reference's long double: the distance between its results and
    restated()'s is the results' own sensitivity to intermediate precision."""
    if "orc64" not in _LIBS:
        if not os.path.exists(FP64_PATH):
            raise RuntimeError(f"oracle library missing: {FP64_PATH} (run make -C oracle)")
        _LIBS["orc64"] = _Lib(FP64_PATH, "orc")
    return _LIBS["orc64"]


def reference_available() -> bool:
    return os.path.exists(REF_PATH)


def reference() -> "_Lib":
    if "ref" not in _LIBS:
        if not os.path.exists(REF_PATH):
            raise RuntimeError(f"reference build missing: {REF_PATH} (run make -C oracle ref)")
        _LIBS["ref"] = _Lib(REF_PATH, "ref")
    return _LIBS["ref"]


def material(m) -> Material:
    return Material(*[float(x) for x in m.astuple()])


class PhaseOracle:
    """Scalar / batch eutectic evaluation through one of the two libraries."""

    def __init__(self, mat, lib: _Lib | None = None):
        self.lib = lib or restated()
        self.mat = material(mat)

    def derived(self) -> dict:
        d = Derived()
        code = self.lib.f("phase_derive")(C.byref(self.mat), C.byref(d))
        if code:
            raise ValueError(f"invalid material parameters (class {code})")
        return {n: getattr(d, n) for n, _ in Derived._fields_}

    def boundaries(self, Cc: float, P: float):
        b = Bounds()
        code = self.lib.f("phase_boundaries")(C.byref(self.mat), C.c_double(Cc), C.c_double(P), C.byref(b))
        return code, {n: getattr(b, n) for n, _ in Bounds._fields_}

    def evaluate(self, H: float, Cc: float, P: float):
        s = Phase()
        code = self.lib.f("phase_evaluate")(C.byref(self.mat), C.c_double(H), C.c_double(Cc), C.c_double(P), C.byref(s))
        return code, {n: getattr(s, n) for n, _ in Phase._fields_}

    def classify(self, H: float, Cc: float, P: float):
        r = C.c_int(0)
        code = self.lib.f("phase_classify")(C.byref(self.mat), C.c_double(H), C.c_double(Cc), C.c_double(P), C.byref(r))
        return code, r.value

    def evaluate_batch(self, H, Cc, P=None, P_const=0.0):
        H = np.ascontiguousarray(H, dtype=np.float64)
        Cc = np.ascontiguousarray(Cc, dtype=np.float64)
        P = None if P is None else np.ascontiguousarray(P, dtype=np.float64)
        out = np.zeros(H.size, dtype=PHASE_DTYPE)
        bad = C.c_longlong(-1)
        code = self.lib.f("phase_evaluate_batch")(
            C.byref(self.mat), _dptr(H), _dptr(Cc), _dptr(P), C.c_double(P_const), C.c_size_t(H.size),
            out.ctypes.data_as(C.c_void_p), C.byref(bad))
        return code, bad.value, out


def transport_opts(w, *, uniform_tables=False, threads=0, integrator=None, pressure=0.0,
                   dt_initial=1e30, dt_max=1e30, dt_min=1e-14, cfl=None, inflow_H=1.0, H_policy=0,
                   inflow_C=0.3, C_policy=0, lf_global=0, lf_global_speed=0.0, mesh_family=0, perturbation=0.0,
                   mesh_seed=1, theta=0.0) -> TransportOpts:
    return TransportOpts(nx=w.nx, ny=w.ny, x0=w.x0, x1=w.x1, y0=w.y0, y1=w.y1, pressure=pressure,
                         cfl=w.cfl if cfl is None else cfl, dt_initial=dt_initial, dt_max=dt_max,
                         dt_min=dt_min, theta=float(theta), inflow_H=inflow_H, inflow_C=inflow_C, H_policy=int(H_policy),
                         C_policy=int(C_policy), integrator=int(integrator if integrator is not None else w.integrator),
                         lf_global=int(lf_global), lf_global_speed=float(lf_global_speed),
                         uniform_tables=int(uniform_tables), threads=int(threads),
                         mesh_family=int(mesh_family), perturbation=float(perturbation), seed=int(mesh_seed))


class TransportOracle:
    """One transport instance of the CPU oracle (restated or reference-backed)."""

    def __init__(self, mat, w, lib: _Lib | None = None, **kw):
        self.lib = lib or restated()
        self.w = w
        self.mat = material(mat)
        self.opts = transport_opts(w, **kw)
        self.h = self.lib.f("transport_create")(C.byref(self.mat), C.byref(self.opts))
        if not self.h:
            raise RuntimeError("oracle transport setup failed")

    def close(self):
        if self.h:
            self.lib.f("transport_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_face_velocity(self, vs, ud):
        self._vs = np.ascontiguousarray(vs, dtype=np.float64)
        self._ud = np.ascontiguousarray(ud, dtype=np.float64)
        return self.lib.f("transport_set_face_velocity")(self.h, _dptr(self._vs), _dptr(self._ud))

    def set_state(self, H, Cc, time=0.0):
        H = np.ascontiguousarray(H, dtype=np.float64)
        Cc = np.ascontiguousarray(Cc, dtype=np.float64)
        return self.lib.f("transport_set_state")(self.h, _dptr(H), _dptr(Cc), C.c_double(time))

    def get_state(self):
        n = self.w.cells
        H, Cc, T, phi = (np.zeros(n) for _ in range(4))
        self.lib.f("transport_get_state")(self.h, _dptr(H), _dptr(Cc), _dptr(T), _dptr(phi))
        return H, Cc, T, phi

    def rhs(self):
        n = self.w.cells
        rh, rc, T, phi, rate = (np.zeros(n) for _ in range(5))
        rep = StepReport()
        code = self.lib.f("transport_rhs")(self.h, _dptr(rh), _dptr(rc), _dptr(T), _dptr(phi), _dptr(rate), C.byref(rep))
        return code, dict(rhsH=rh, rhsC=rc, T=T, phi=phi, rate=rate,
                          **{n: getattr(rep, n) for n, _ in StepReport._fields_})

    def limiter(self):
        n = self.w.cells
        a, b = np.zeros(n), np.zeros(n)
        code = self.lib.f("transport_limiter")(self.h, _dptr(a), _dptr(b))
        return code, a, b

    def set_diffusion(self, kappa: float, types=(0, 0, 0, 0), values=(0.0, 0.0, 0.0, 0.0)):
        """kappa and per-wall thermal conditions (bottom, top, left, right):
        0 zero flux, 1 prescribed temperature, 2 prescribed outward flux."""
        ti = (C.c_int * 4)(*[int(x) for x in types])
        tv = (C.c_double * 4)(*[float(x) for x in values])
        return self.lib.f("transport_set_diffusion")(self.h, float(kappa), ti, tv)

    def set_pressure_model(self, model: int, value: float):
        """0: constant pressure `value` Pa; 1: lithostatic with the surface at y = value."""
        return self.lib.f("transport_set_pressure_model")(self.h, int(model), float(value))

    def set_cell_velocity(self, vs_y, ud_y):
        a = np.ascontiguousarray(vs_y, dtype=np.float64)
        b = np.ascontiguousarray(ud_y, dtype=np.float64)
        self._cellv = (a, b)
        return self.lib.f("transport_set_cell_velocity")(self.h, _dptr(a), _dptr(b))

    def vertices(self) -> np.ndarray:
        xy = np.zeros(2 * (self.w.nx + 1) * (self.w.ny + 1))
        self.lib.f("transport_vertices")(self.h, _dptr(xy))
        return xy

    def set_time_control(self, control: int, t_end: float = float("inf")):
        return self.lib.f("transport_set_time_control")(self.h, int(control), float(t_end))

    def step(self, nsteps: int):
        reps = (StepReport * max(1, nsteps))()
        code = self.lib.f("transport_step")(self.h, C.c_int(nsteps), reps)
        return code, [{n: getattr(r, n) for n, _ in StepReport._fields_} for r in reps[:nsteps]]

    # Legacy dry preheat (src/couple/preheat.cpp) on this instance: velocity =
    # vs of set_face_velocity, kappa and walls of set_diffusion, control and
    # time.end of set_time_control.
    def preheat_begin(self):
        rate = np.zeros(self.w.cells)
        limit = C.c_double()
        first = PreheatStep()
        code = self.lib.f("preheat_begin")(self.h, _dptr(rate), C.byref(limit), C.byref(first))
        return code, rate, limit.value, _row(first)

    def preheat_rhs(self):
        rhs = np.zeros(self.w.cells)
        b = C.c_double()
        code = self.lib.f("preheat_rhs")(self.h, _dptr(rhs), C.byref(b))
        return code, rhs, b.value

    def preheat_advance(self, nsteps: int, max_steps: int = 1 << 62):
        rows = (PreheatStep * max(1, nsteps))()
        taken = C.c_longlong()
        code = self.lib.f("preheat_advance")(self.h, C.c_longlong(max_steps), C.c_longlong(nsteps), rows,
                                             C.byref(taken))
        return code, [_row(r) for r in rows[:taken.value]]

    def preheat_diagnostics(self):
        T, phi = np.zeros(self.w.cells), np.zeros(self.w.cells)
        code = self.lib.f("preheat_diagnostics")(self.h, _dptr(T), _dptr(phi))
        return code, T, phi

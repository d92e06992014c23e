"""ctypes binding of the mantlepar_b200 C ABI (include/mantlepar/mp.h).

The CUDA library is loaded from the package directory; there is no CPU
fallback: if it is missing, importing the bindings fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# MP_CHECKED=1 loads the bounds-checked build (python -m mantlepar_b200.build --checked).
LIB_PATH = os.path.join(HERE, "libmantlepar_b200_checked.so" if os.environ.get("MP_CHECKED") == "1"
                        else "libmantlepar_b200.so")
HEADER = os.path.join(ROOT, "include", "mantlepar", "mp.h")

STATUS = {
    0: "MP_OK", 60: "MP_ERR_ARG_SIZ", 62: "MP_ERR_ARG_WRONG", 63: "MP_ERR_ARG_OUTOFRANGE",
    72: "MP_ERR_FP", 73: "MP_ERR_ARG_WRONGSTATE", 77: "MP_ERR_PLIB", 91: "MP_ERR_NOT_CONVERGED",
    101: "MP_ERR_PHASE_INVALID", 102: "MP_ERR_PHASE_OVERFLOW", 103: "MP_ERR_PHASE_RUNTIME",
    110: "MP_ERR_TIMEOUT", 111: "MP_ERR_NOMEM", 112: "MP_ERR_CUDA",
}


class MPError(RuntimeError):
    """A failed mantlepar_b200 call; `code` is the mp_status value."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


class Material(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ["Tm0", "Te0", "nu", "L", "cp", "Xe", "rho", "rhor", "mus", "mul", "k0", "g", "alpha0"]]


class Derived(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ["dT", "h0", "gamma", "LD", "TDm0", "TDe0", "invk0", "l0", "u0", "p0", "t0"]]


class Bounds(C.Structure):
    _fields_ = [(n, C.c_double) for n in ["Tep", "Tmp", "H_eutectic_end", "H_liquidus"]]


class PhaseSoA(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in
                ["phi1", "phi2", "phil", "cl", "cs", "TDp", "Tep", "dTD_dCD", "dTD_dHD", "region", "flags"]]


class MeshDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("x0", C.c_double), ("x1", C.c_double),
                ("y0", C.c_double), ("y1", C.c_double)]


class TransportOpts(C.Structure):
    _fields_ = [("material", Material), ("pressure", C.c_double), ("cfl", C.c_double),
                ("dt_initial", C.c_double), ("dt_max", C.c_double), ("dt_min", C.c_double),
                ("theta", C.c_double), ("inflow_H", C.c_double), ("inflow_C", C.c_double),
                ("H_policy", C.c_int), ("C_policy", C.c_int), ("integrator", C.c_int),
                ("lf_global", C.c_int), ("lf_global_speed", C.c_double), ("diffusivity", C.c_double),
                ("precision", C.c_int)]


class StepReport(C.Structure):
    _fields_ = [("status", C.c_int), ("retries", C.c_int), ("dt", C.c_double), ("time", C.c_double),
                ("courant", C.c_double), ("boundaryH", C.c_double), ("boundaryC", C.c_double),
                ("sourceH", C.c_double), ("maxRate", C.c_double), ("divergence", C.c_double),
                ("balanceH", C.c_double), ("balanceC", C.c_double), ("H_integral", C.c_double),
                ("C_integral", C.c_double)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("accepted", C.c_int), ("time", C.c_double), ("queue_s", C.c_double),
                ("latency_s", C.c_double), ("cells", C.c_double)]


class StageTotals(C.Structure):
    _fields_ = [(n, C.c_double) for n in ["boundaryH", "boundaryC", "sourceH", "maxRate", "divergence"]]


class PreheatOpts(C.Structure):
    _fields_ = [("material", Material), ("pressure_model", C.c_int), ("pressure", C.c_double),
                ("end", C.c_double), ("max_steps", C.c_longlong), ("control", C.c_int),
                ("dt_initial", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double), ("cfl", C.c_double),
                ("diffusivity", C.c_double), ("thermal_type", C.c_int * 4), ("thermal_value", C.c_double * 4),
                ("H_policy", C.c_int), ("inflow_H", C.c_double), ("lf_global", C.c_int),
                ("lf_global_speed", C.c_double)]


class PreheatStep(C.Structure):
    _fields_ = [("step", C.c_longlong), ("time", C.c_double), ("dt", C.c_double), ("courant", C.c_double),
                ("integral", C.c_double), ("minimum", C.c_double), ("maximum", C.c_double),
                ("boundaryFlux", C.c_double), ("balanceError", C.c_double)]


class PreheatReport(C.Structure):
    _fields_ = [(n, C.c_double) for n in ["initialTime", "finalTime", "stepLimit", "initialIntegral",
                                          "finalIntegral", "boundaryIntegral"]]


_lib = None


def lib() -> C.CDLL:
    """Load (once) the CUDA library; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"mantlepar_b200 CUDA library missing: {LIB_PATH} "
                           "(build it with `python -m mantlepar_b200.build`)")
    L = C.CDLL(LIB_PATH)
    vp, dp, i, d, sz = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_double, C.c_size_t
    sig = {
        "mp_last_error_string": (C.c_char_p, []),
        "mp_kernel_launches": (C.c_ulonglong, []),
        "mp_phase_create": (i, [C.POINTER(Material), C.POINTER(vp)]),
        "mp_phase_set_params": (i, [vp, C.POINTER(Material)]),
        "mp_phase_get_params": (i, [vp, C.POINTER(Material)]),
        "mp_phase_get_derived": (i, [vp, C.POINTER(Derived)]),
        "mp_phase_destroy": (None, [vp]),
        "mp_phase_boundaries": (i, [vp, d, d, C.POINTER(Bounds)]),
        "mp_phase_evaluate_batch": (i, [vp, vp, vp, vp, d, sz, C.POINTER(PhaseSoA), C.POINTER(C.c_longlong), vp]),
        "mp_phase_evaluate_host": (i, [vp, vp, vp, vp, d, sz, C.POINTER(PhaseSoA), C.POINTER(C.c_longlong)]),
        "mp_phase_pressure_corrected_temperature": (i, [vp, d, d, dp]),
        "mp_phase_static_pressure": (i, [vp, d, d, dp]),
        "mp_transport_create": (i, [C.POINTER(MeshDesc), C.POINTER(TransportOpts), vp, C.POINTER(vp)]),
        "mp_transport_destroy": (None, [vp]),
        "mp_transport_set_face_velocity": (i, [vp, vp, vp]),
        "mp_transport_set_state": (i, [vp, vp, vp, d]),
        "mp_transport_get_state": (i, [vp, vp, vp, vp, vp]),
        "mp_transport_rhs": (i, [vp, vp, vp, vp, vp, vp, C.POINTER(StageTotals)]),
        "mp_transport_step": (i, [vp, i, C.POINTER(StepReport)]),
        "mp_transport_limiter": (i, [vp, vp, vp]),
        "mp_transport_set_device_steps": (i, [vp, i]),
        "mp_transport_run_stats": (i, [vp, C.POINTER(C.c_ulonglong)]),
        "mp_batch_set_device_steps": (i, [vp, i]),
        "mp_batch_set_cell_velocity": (i, [vp, i, vp, vp]),
        "mp_batch_run_stats": (i, [vp, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
        "mp_transport_profile": (i, [vp, i]),
        "mp_transport_kernel_times": (i, [vp, C.POINTER(C.c_double), C.POINTER(C.c_ulonglong)]),
        "mp_probe_fp64_peak": (i, [vp, C.POINTER(C.c_double)]),
        "mp_transport_rhs_noalloc": (i, [C.POINTER(MeshDesc), C.POINTER(TransportOpts), vp, vp, vp, vp,
                                         vp, vp, vp, vp, vp, C.POINTER(StageTotals), vp]),
        "mp_batch_create": (i, [C.POINTER(MeshDesc), i, C.POINTER(TransportOpts), vp, C.POINTER(vp)]),
        "mp_batch_destroy": (None, [vp]),
        "mp_batch_add": (i, [vp, C.POINTER(MeshDesc), C.POINTER(C.c_int)]),
        "mp_batch_remove": (i, [vp, i]),
        "mp_batch_instance_bytes": (sz, [C.POINTER(MeshDesc)]),
        "mp_batch_add_quads": (i, [vp, C.POINTER(MeshDesc), vp, C.POINTER(i)]),
        "mp_batch_bytes_in_use": (sz, [vp]),
        "mp_batch_slots": (i, [vp]),
        "mp_batch_set_face_velocity": (i, [vp, i, vp, vp]),
        "mp_batch_set_state": (i, [vp, i, vp, vp, d]),
        "mp_batch_get_state": (i, [vp, i, vp, vp, vp, vp, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "mp_batch_step": (i, [vp, i, C.POINTER(StepReport)]),
        "mp_batch_autotune": (i, [vp, i, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        "mp_batch_profile": (i, [vp, i]),
        "mp_batch_set_end_time": (i, [vp, i, d]),
        "mp_batch_finished": (i, [vp, i]),
        "mp_serve_create": (i, [C.POINTER(TransportOpts), sz, C.POINTER(vp)]),
        "mp_serve_destroy": (None, [vp]),
        "mp_serve_submit": (i, [vp, C.POINTER(MeshDesc), vp, vp, vp, vp, d, C.POINTER(C.c_longlong)]),
        "mp_serve_submit_quads": (i, [vp, C.POINTER(MeshDesc), vp, vp, vp, vp, vp, d, C.POINTER(C.c_longlong)]),
        "mp_serve_wait": (i, [vp, C.c_longlong, d, vp, vp, vp, vp, C.POINTER(RequestInfo)]),
        "mp_serve_stats": (i, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                               C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "mp_serve_set_policy": (i, [vp, i, d]),
        "mp_transport_set_time_control": (i, [vp, i, d]),
        "mp_transport_set_thermal_bc": (i, [vp, C.POINTER(C.c_int), dp]),
        "mp_transport_set_pressure_model": (i, [vp, i, d]),
        "mp_transport_set_cell_velocity": (i, [vp, vp, vp]),
        "mp_batch_set_thermal_bc": (i, [vp, C.POINTER(C.c_int), dp]),
        "mp_transport_create_slab": (i, [C.POINTER(MeshDesc), i, i, C.POINTER(TransportOpts), vp, C.POINTER(vp)]),
        "mp_transport_slab_layout": (i, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]),
        "mp_transport_set_hooks": (i, [vp, vp, vp, vp]),
        "mp_transport_get_time": (i, [vp, dp, C.POINTER(C.c_int)]),
        "mp_batch_kernel_times": (i, [vp, C.POINTER(C.c_double), C.POINTER(C.c_ulonglong)]),
        "mp_transport_create_quads": (i, [C.POINTER(MeshDesc), vp, C.POINTER(TransportOpts), vp, C.POINTER(vp)]),
        "mp_transport_instance_bytes": (sz, [C.POINTER(MeshDesc), i]),
        "mp_mesh_vertices": (i, [C.POINTER(MeshDesc), i, d, C.c_ulonglong, vp]),
        "mp_transport_create_quads_slab": (i, [C.POINTER(MeshDesc), vp, i, i, C.POINTER(TransportOpts), vp,
                                               C.POINTER(vp)]),
        "mp_preheat_create": (i, [C.POINTER(MeshDesc), C.POINTER(PreheatOpts), vp, C.POINTER(vp)]),
        "mp_preheat_create_quads": (i, [C.POINTER(MeshDesc), vp, C.POINTER(PreheatOpts), vp, C.POINTER(vp)]),
        "mp_preheat_destroy": (None, [vp]),
        "mp_preheat_set_velocity": (i, [vp, vp]),
        "mp_preheat_set_state": (i, [vp, vp, vp, d, C.c_longlong]),
        "mp_preheat_get_state": (i, [vp, vp, dp, C.POINTER(C.c_longlong)]),
        "mp_preheat_begin": (i, [vp, vp, dp, C.POINTER(PreheatStep)]),
        "mp_preheat_rhs": (i, [vp, vp, dp]),
        "mp_preheat_advance": (i, [vp, C.c_longlong, C.POINTER(PreheatStep), C.POINTER(C.c_longlong)]),
        "mp_preheat_diagnostics": (i, [vp, vp, vp]),
        "mp_preheat_run": (i, [vp, C.POINTER(PreheatReport), C.POINTER(PreheatStep), C.c_longlong,
                               C.POINTER(C.c_longlong), vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(code: int) -> None:
    if code != 0:
        raise MPError(code, lib().mp_last_error_string().decode())


def header_functions() -> list[str]:
    """Names of the functions declared in include/mantlepar/mp.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mp_[a-z0-9_]+)\s*\(", text)))


def kernel_launches() -> int:
    return int(lib().mp_kernel_launches())

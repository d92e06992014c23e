"""Host mirror of mantle::phase::EutecticModel over the CUDA phase kernel.

Same names, argument meaning and error behaviour as
src/phase/eutectic_rescaled.h:103-136: invalid input raises ValueError
(std::invalid_argument), unrepresentable scales/temperatures OverflowError
(std::overflow_error), fractions outside [0,1] RuntimeError
(std::runtime_error); a rejected setParameters leaves the model unchanged.
Evaluation always runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np
import torch

from . import _capi
from .synthetic import Material as MaterialParameters

FIELDS = ["phi1", "phi2", "phil", "cl", "cs", "TDp", "Tep", "dTD_dCD", "dTD_dHD"]
REGIONS = {1: "PureSolid", 2: "TwoSolids", 3: "Eutectic", 4: "SolidLiquid", 5: "Liquid", 6: "PureMelting"}


@dataclasses.dataclass
class PhaseState:
    phi1: float = 0.0
    phi2: float = 0.0
    phil: float = 0.0
    cl: float = 0.0
    cs: float = 0.0
    region: int = 1
    TDp: float = 0.0
    Tep: float = 0.0
    dTD_dCD: float = 0.0
    dTD_dHD: float = 0.0
    has_solid: bool = False
    has_liquid: bool = False
    finite_temperature_derivatives: bool = True


@dataclasses.dataclass
class PhaseBoundaries:
    Tep: float
    Tmp: float
    H_eutectic_end: float
    H_liquidus: float


def _raise(code: int) -> None:
    if code == 0:
        return
    msg = _capi.lib().mp_last_error_string().decode()
    if code == 101:
        raise ValueError(msg)
    if code == 102:
        raise OverflowError(msg)
    if code == 103:
        raise RuntimeError(msg)
    raise _capi.MPError(code, msg)


def _material(p: MaterialParameters) -> _capi.Material:
    return _capi.Material(*[float(x) for x in dataclasses.astuple(p)])


class EutecticModel:
    """Binary eutectic equilibrium (component-1-rich side, 0 <= CD <= Xe)."""

    def __init__(self, parameters: MaterialParameters | None = None, device: int | None = None):
        self._lib = _capi.lib()
        self._device = torch.device("cuda", device if device is not None else torch.cuda.current_device())
        p = parameters if parameters is not None else MaterialParameters()
        h = C.c_void_p()
        m = _material(p)
        _raise(self._lib.mp_phase_create(C.byref(m), C.byref(h)))
        self._h = h
        self._params = dataclasses.replace(p)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.mp_phase_destroy(h)
            self._h = None

    def parameters(self) -> MaterialParameters:
        return dataclasses.replace(self._params)

    def derived(self) -> dict:
        d = _capi.Derived()
        _raise(self._lib.mp_phase_get_derived(self._h, C.byref(d)))
        return {n: getattr(d, n) for n, _ in _capi.Derived._fields_}

    def setParameters(self, p: MaterialParameters) -> None:
        m = _material(p)
        _raise(self._lib.mp_phase_set_params(self._h, C.byref(m)))
        self._params = dataclasses.replace(p)

    set_parameters = setParameters

    def boundaries(self, CD: float, P: float) -> PhaseBoundaries:
        b = _capi.Bounds()
        _raise(self._lib.mp_phase_boundaries(self._h, float(CD), float(P), C.byref(b)))
        return PhaseBoundaries(b.Tep, b.Tmp, b.H_eutectic_end, b.H_liquidus)

    def evaluate_batch(self, H, Cc, P=None, P_const: float = 0.0, fields=None, raise_on_error: bool = True):
        """Evaluate many points on the GPU.

        H, Cc (and P) are array-likes or CUDA tensors of equal length. Returns
        (outputs, status, first_bad); outputs maps each requested field name
        (FIELDS + "region" + "flags") to a CUDA tensor.
        """
        dev = self._device
        Ht = torch.as_tensor(H, dtype=torch.float64, device=dev).contiguous()
        Ct = torch.as_tensor(Cc, dtype=torch.float64, device=dev).contiguous()
        Pt = None if P is None else torch.as_tensor(P, dtype=torch.float64, device=dev).contiguous()
        n = Ht.numel()
        want = fields if fields is not None else FIELDS + ["region", "flags"]
        out = {}
        soa = _capi.PhaseSoA()
        for f in want:
            if f == "region":
                t = torch.empty(n, dtype=torch.int8, device=dev)
            elif f == "flags":
                t = torch.empty(n, dtype=torch.uint8, device=dev)
            else:
                t = torch.empty(n, dtype=torch.float64, device=dev)
            out[f] = t
            setattr(soa, f, t.data_ptr())
        bad = C.c_longlong(-1)
        stream = torch.cuda.current_stream(dev).cuda_stream
        code = self._lib.mp_phase_evaluate_batch(
            self._h, Ht.data_ptr(), Ct.data_ptr(), Pt.data_ptr() if Pt is not None else None,
            float(P_const), n, C.byref(soa), C.byref(bad), stream)
        if raise_on_error:
            _raise(code)
        return out, code, bad.value

    def evaluate(self, HD: float, CD: float, P: float) -> PhaseState:
        out, _, _ = self.evaluate_batch(np.array([HD]), np.array([CD]), np.array([P]))
        v = {k: out[k].cpu().numpy()[0] for k in out}
        flags = int(v["flags"])
        return PhaseState(phi1=float(v["phi1"]), phi2=float(v["phi2"]), phil=float(v["phil"]), cl=float(v["cl"]),
                          cs=float(v["cs"]), region=int(v["region"]), TDp=float(v["TDp"]), Tep=float(v["Tep"]),
                          dTD_dCD=float(v["dTD_dCD"]), dTD_dHD=float(v["dTD_dHD"]), has_solid=bool(flags & 1),
                          has_liquid=bool(flags & 2), finite_temperature_derivatives=bool(flags & 4))

    def classify(self, HD: float, CD: float, P: float) -> int:
        """Region only (eutectic_rescaled.cpp:187-190): a failure of the
        evaluation after the region was selected still returns the region."""
        out, code, _ = self.evaluate_batch(np.array([HD]), np.array([CD]), np.array([P]), fields=["region"],
                                           raise_on_error=False)
        region = int(out["region"].cpu().numpy()[0])
        if code and not (region and code in (102, 103)):
            _raise(code)
        return region

    def pressureCorrectedTemperature(self, TD: float, P: float) -> float:
        v = C.c_double(0.0)
        _raise(self._lib.mp_phase_pressure_corrected_temperature(self._h, float(TD), float(P), C.byref(v)))
        return v.value

    def staticPressure(self, zD: float, length_scale: float | None = None) -> float:
        ls = self.derived()["l0"] if length_scale is None else float(length_scale)
        v = C.c_double(0.0)
        _raise(self._lib.mp_phase_static_pressure(self._h, float(zD), ls, C.byref(v)))
        return v.value

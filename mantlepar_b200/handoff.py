"""Handoff files of the coupled transport, as the reference writes and reads them.

* `cellH1.dat` / `cellC1.dat`: cell averages in natural order j*nx + i, one
  mesh row per line, values separated by one space, 17 significant digits
  (src/couple/initialization.cpp:645-680);
* `transport_state.json`: the manifest that describes them (schema 1,
  initialization.cpp:823-840) and that LoadPreheatState checks before it
  imports a state (src/couple/evolve.cpp:54-125);
* `evolution_history.csv`: one row per accepted step with the reference's
  columns (evolve.cpp:443, WriteRow :399-426).

Files are written to a temporary name and renamed, so a reader never sees a
partial file. The names, keys, units strings and validation rules are the
reference's, so a state can pass between this library and a reference run.
"""
from __future__ import annotations

import dataclasses
import json
import math
import os

import numpy as np

HISTORY_COLUMNS = ("step,time,time_years,dt,courant,H_integral,C_integral,h_mean_J_kg,C_mean,h_min_J_kg,"
                   "h_max_J_kg,C_min,C_max,phi_min,phi_max,outward_H_flux,outward_C_flux,adiabatic_H_source,"
                   "H_balance_error,C_balance_error,mixture_divergence_max,flow_relative_residual,retries")
SECONDS_PER_YEAR = 365 * 24 * 3600


class HandoffError(ValueError):
    """A handoff file is missing, malformed or does not match the run."""


@dataclasses.dataclass
class MeshInfo:
    nx: int
    ny: int
    domain: tuple[float, float, float, float]      # x0, x1, y0, y1
    family: str = "rectangular"
    perturbation: float = 0.0
    seed: int = 0

    @classmethod
    def of(cls, w) -> "MeshInfo":
        return cls(w.nx, w.ny, (w.x0, w.x1, w.y0, w.y1))


def _g17(v: float) -> str:
    return format(float(v), ".17g")


def _atomic_write(path: str, text: str) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write(text)
    os.replace(tmp, path)


def _matrix_text(a: np.ndarray, nx: int) -> str:
    rows = np.asarray(a, dtype=np.float64).reshape(-1, nx)
    return "".join(" ".join(_g17(v) for v in row) + "\n" for row in rows)


def write_state(directory: str, mesh: MeshInfo, H, C, time: float, accepted_steps: int, derived: dict) -> None:
    """cellH1.dat, cellC1.dat and transport_state.json of a state."""
    n = mesh.nx * mesh.ny
    H, C = np.asarray(H, dtype=np.float64).ravel(), np.asarray(C, dtype=np.float64).ravel()
    if H.size != n or C.size != n:
        raise HandoffError(f"fields hold {H.size}/{C.size} values, the mesh has {n} cells")
    os.makedirs(directory, exist_ok=True)
    _atomic_write(os.path.join(directory, "cellH1.dat"), _matrix_text(H, mesh.nx))
    _atomic_write(os.path.join(directory, "cellC1.dat"), _matrix_text(C, mesh.nx))
    manifest = {
        "schema_version": 1, "status": "complete",
        "representation": "cell averages", "ordering": "j*nx+i",
        "H": {"file": "cellH1.dat", "units": "h/(cp*dT)"},
        "C": {"file": "cellC1.dat", "units": "fraction"},
        "time": float(time), "time_s": float(time) * derived["t0"],
        "accepted_steps": int(accepted_steps),
        "mesh": {"family": mesh.family, "nx": mesh.nx, "ny": mesh.ny, "domain": [float(x) for x in mesh.domain],
                 "perturbation": float(mesh.perturbation), "seed": int(mesh.seed)},
        "scales": {"enthalpy_Jkg": derived["h0"], "length_m": derived["l0"], "time_s": derived["t0"]},
    }
    _atomic_write(os.path.join(directory, "transport_state.json"), json.dumps(manifest, indent=1) + "\n")


def _require(ok: bool, msg: str) -> None:
    if not ok:
        raise HandoffError(msg)


def _close(a: float, b: float) -> bool:
    return math.isfinite(a) and abs(a - b) <= 1e-12 * max(1.0, abs(a), abs(b))


def read_state(directory: str, mesh: MeshInfo, derived: dict, Xe: float):
    """Validate and import a state as LoadPreheatState does (evolve.cpp:54-125).

    Returns (H, C, source_time)."""
    path = os.path.join(directory, "transport_state.json")
    try:
        with open(path) as f:
            m = json.load(f)
    except (OSError, ValueError) as e:
        raise HandoffError(f"cannot read {path}: {e}") from e
    try:
        _require(m["schema_version"] == 1 and m["status"] == "complete", "Preheat manifest must be complete schema 1")
        _require(m["representation"] == "cell averages" and m["ordering"] == "j*nx+i",
                 "Unsupported preheat representation/order")
        _require(m["H"]["units"] == "h/(cp*dT)" and m["C"]["units"] == "fraction", "Preheat units do not match")
        _require(m["H"]["file"] == "cellH1.dat" and m["C"]["file"] == "cellC1.dat", "Unsupported preheat filenames")
        mm = m["mesh"]
        _require(mm["family"] == mesh.family and int(mm["nx"]) == mesh.nx and int(mm["ny"]) == mesh.ny,
                 "Preheat mesh does not match evolution mesh")
        for k in range(4):
            _require(_close(float(mm["domain"][k]), mesh.domain[k]), "Preheat domain does not match")
        if mesh.family != "rectangular":
            _require(_close(float(mm["perturbation"]), mesh.perturbation) and int(mm["seed"]) == mesh.seed,
                     "Preheat mesh perturbation does not match")
        sc = m["scales"]
        _require(_close(float(sc["enthalpy_Jkg"]), derived["h0"]) and _close(float(sc["length_m"]), derived["l0"])
                 and _close(float(sc["time_s"]), derived["t0"]),
                 "Preheat scales do not match; explicit physical conversion is required")
        source_time = float(m["time"])
        _require(math.isfinite(source_time), "Nonfinite source time")
    except (KeyError, TypeError, ValueError) as e:
        if isinstance(e, HandoffError):
            raise
        raise HandoffError(f"malformed preheat manifest: {e}") from e
    n = mesh.nx * mesh.ny
    out = []
    for k, name in enumerate(("cellH1.dat", "cellC1.dat")):
        try:
            with open(os.path.join(directory, name)) as f:
                tokens = f.read().split()
        except OSError as e:
            raise HandoffError("Cannot open preheat field") from e
        _require(len(tokens) >= n, "Incomplete preheat cell-average matrix")
        _require(len(tokens) == n, "Extra entries in preheat cell-average matrix")
        try:
            v = np.array([float(t) for t in tokens])
        except ValueError as e:
            raise HandoffError("Incomplete preheat cell-average matrix") from e
        _require(bool(np.all(np.isfinite(v)) and np.all(v >= 0) and (k == 0 or np.all(v <= Xe))),
                 "Inadmissible preheat cell average")
        out.append(v)
    return out[0], out[1], source_time


class HistoryWriter:
    """evolution_history.csv rows (WriteRow, evolve.cpp:399-426)."""

    def __init__(self, path: str, mesh: MeshInfo, derived: dict):
        self.f = open(path, "w")
        self.f.write(HISTORY_COLUMNS + "\n")
        self.f.flush()
        self.mesh, self.d = mesh, derived
        x0, x1, y0, y1 = mesh.domain
        self.area = (x1 - x0) * (y1 - y0)
        self.cell_area = self.area / (mesh.nx * mesh.ny)

    def row(self, step: int, time: float, H, C, phi, report: dict | None = None, dt: float = 0.0,
            courant: float = 0.0, retries: int = 0, flow_residual: float = 0.0) -> None:
        """One accepted state: report holds the step report's boundary fluxes,
        source, balance errors and divergence (zeros for the initial row)."""
        r = report or {}
        H, C, phi = (np.asarray(a, dtype=np.float64) for a in (H, C, phi))
        Hi, Ci = float(np.sum(H * self.cell_area)), float(np.sum(C * self.cell_area))
        d = self.d
        vals = [time, time * d["t0"] / SECONDS_PER_YEAR, dt, courant, Hi, Ci, Hi / self.area * d["h0"],
                Ci / self.area, H.min() * d["h0"], H.max() * d["h0"], C.min(), C.max(), phi.min(), phi.max(),
                r.get("boundaryH", 0.0), r.get("boundaryC", 0.0), r.get("sourceH", 0.0), r.get("balanceH", 0.0),
                r.get("balanceC", 0.0), r.get("divergence", 0.0), flow_residual]
        self.f.write(f"{int(step)}," + ",".join(_g17(v) for v in vals) + f",{int(retries)}\n")
        self.f.flush()

    def close(self):
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def read_history(path: str) -> list[dict]:
    with open(path) as f:
        header = f.readline().strip()
        _require(header == HISTORY_COLUMNS, "unexpected evolution_history.csv header")
        cols = header.split(",")
        rows = []
        for line in f:
            parts = line.strip().split(",")
            rows.append({c: (int(p) if c in ("step", "retries") else float(p)) for c, p in zip(cols, parts)})
    return rows

"""Generate the committed golden fixtures from the REFERENCE's own code.

Run in a container where the reference sources are mounted (they are not on
GPU machines):

    make -C oracle ref            # compiles the reference's sources into oracle/_ref
    python tests/golden/make_golden.py [phase] [transport] [preheat] [quads]

Writes, next to this script:
  phase_golden.npz      inputs and EutecticModel::evaluate outputs of the
                        reference (src/phase/eutectic_rescaled.cpp) for the
                        three parameter sets x four pressures of its own test:
                        interval-end nextafter neighbours, forward-constructed
                        known answers, seeded random states, invalid inputs.
  transport_golden.npz  the reference-backed transport oracle (the reference's
                        Reconstruction/TensorStencilPoly/diffusion sampling/
                        EutecticModel under the restated evolve.cpp driver) on
                        seeded synthetic workloads: one RHS and short runs on
                        20x20 and on small meshes with every boundary class,
                        plus 200-step SSPRK2 and SSPRK3 runs of 20x20.
  preheat_golden.npz    the reference-backed legacy dry preheat on the seeded
                        cases of tests/preheat_cases.py.
  quads_golden.npz      the reference-backed transport on perturbed-quadrilateral
                        and sine-stretched meshes: RHS, limiter, 10 SSPRK3 steps.
Arguments (phase, transport, preheat, quads) select fixtures; none = all.
"""
from __future__ import annotations

import dataclasses
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import pyoracle as po  # noqa: E402
from mantlepar_b200 import synthetic as sy  # noqa: E402
import phase_known_answers as ka  # noqa: E402


class _RefModel:
    """EutecticModel-shaped view of the reference build (for case generation)."""

    def __init__(self, p):
        self.p = p
        self.o = po.PhaseOracle(p, po.reference())

    def derived(self):
        return self.o.derived()

    def boundaries(self, C, P):
        code, b = self.o.boundaries(C, P)
        assert code == 0
        return type("B", (), b)


def phase_golden():
    rows = []  # (set, H, C, P)
    for si, p in enumerate(ka.parameter_sets()):
        m = _RefModel(p)
        for P in ka.PRESSURES:
            for H, C, _ in ka.region_cases(m, p, P):
                rows.append((si, H, C, P))
            for C, lo, at, hi in ka.boundary_points(m, p, P):
                rows += [(si, lo, C, P), (si, at, C, P), (si, hi, C, P)]
            H, C = ka.conservation_states(p, P, m, 400, seed=13579 + si * 10 + int(abs(P)) % 7)
            rows += [(si, float(h), float(c), P) for h, c in zip(H, C)]
            # invalid inputs: C > Xe, C < 0, non-finite H
            rows += [(si, 1.0, p.Xe * 1.5, P), (si, 1.0, -1e-3, P), (si, float("nan"), 0.1 * p.Xe, P)]
    arr = np.array(rows, dtype=np.float64)
    sets = arr[:, 0].astype(np.int32)
    H, C, P = arr[:, 1], arr[:, 2], arr[:, 3]
    out = {f: np.zeros(len(rows)) for f in ["phi1", "phi2", "phil", "cl", "cs", "TDp", "Tep", "dTD_dCD", "dTD_dHD"]}
    out["region"] = np.zeros(len(rows), np.int32)
    out["flags"] = np.zeros(len(rows), np.int32)
    status = np.zeros(len(rows), np.int32)
    for si, p in enumerate(ka.parameter_sets()):
        o = po.PhaseOracle(p, po.reference())
        idx = np.nonzero(sets == si)[0]
        for k in idx:
            code, s = o.evaluate(H[k], C[k], P[k])
            status[k] = code
            if code == 0:
                for f in out:
                    if f in ("region", "flags"):
                        continue
                    out[f][k] = s[f]
                out["region"][k] = s["region"]
                out["flags"][k] = s["has_solid"] | (s["has_liquid"] << 1) | (s["finite_temperature_derivatives"] << 2)
            else:
                for f in out:
                    if f not in ("region", "flags"):
                        out[f][k] = np.nan
    params = np.array([dataclasses.astuple(p) for p in ka.parameter_sets()])
    np.savez_compressed(os.path.join(HERE, "phase_golden.npz"), set=sets, H=H, C=C, P=P, status=status,
                        params=params, **out)
    print("phase_golden.npz:", len(rows), "states,", int((status != 0).sum()), "rejected")


def transport_golden():
    mat = sy.material_s()
    data = {}
    cases = [("w20", sy.Workload(nx=20, ny=20)), ("w2x2", sy.Workload(nx=2, ny=2)),
             ("w3x5", sy.Workload(nx=3, ny=5, seed=7)), ("w7x4", sy.Workload(nx=7, ny=4, seed=9, noise_H=0.1))]
    for name, w in cases:
        H, C = sy.initial_state(w)
        vs, ud = sy.face_velocity(w)
        t = po.TransportOracle(mat, w, lib=po.reference(), integrator=2)
        t.set_face_velocity(vs, ud)
        t.set_state(H, C)
        code, r = t.rhs()
        assert code == 0, (name, code)
        code, thH, thC = t.limiter()
        assert code == 0
        for k in ["rhsH", "rhsC", "T", "phi", "rate"]:
            data[f"{name}_rhs_{k}"] = r[k]
        data[f"{name}_rhs_totals"] = np.array([r["boundaryH"], r["boundaryC"], r["maxRate"], r["divergence"]])
        data[f"{name}_thetaH"], data[f"{name}_thetaC"] = thH, thC
        for integ in (2, 3):
            t = po.TransportOracle(mat, w, lib=po.reference(), integrator=integ)
            t.set_face_velocity(vs, ud)
            t.set_state(H, C)
            code, reps = t.step(10)
            assert code == 0, (name, integ, code)
            Hs, Cs, T, phi = t.get_state()
            data[f"{name}_rk{integ}_10"] = np.stack([Hs, Cs, T, phi])
            data[f"{name}_rk{integ}_10_dt"] = np.array([r["dt"] for r in reps])
            data[f"{name}_rk{integ}_10_retries"] = np.array([r["retries"] for r in reps])
    w = sy.plain_small()
    H, C = sy.initial_state(w)
    vs, ud = sy.face_velocity(w)
    for integ in (2, 3):
        t = po.TransportOracle(mat, w, lib=po.reference(), integrator=integ)
        t.set_face_velocity(vs, ud)
        t.set_state(H, C)
        code, reps = t.step(200)
        assert code == 0
        Hs, Cs, T, phi = t.get_state()
        data[f"w20_rk{integ}_200"] = np.stack([Hs, Cs, T, phi])
        data[f"w20_rk{integ}_200_dt"] = np.array([r["dt"] for r in reps])
        data[f"w20_rk{integ}_200_retries"] = np.array([r["retries"] for r in reps])
    np.savez_compressed(os.path.join(HERE, "transport_golden.npz"), **data)
    print("transport_golden.npz:", len(data), "arrays")


ROW_FIELDS = ["step", "time", "dt", "courant", "integral", "minimum", "maximum", "boundaryFlux", "balanceError"]


def preheat_golden():
    """The reference-backed preheat (src/couple/preheat.cpp driver over the
    reference's reconstruction, advective and diffusive flux functions) on the
    seeded cases of tests/preheat_cases.py: Build, one RHS, the whole run and
    the diagnostics."""
    import preheat_cases as pc
    data = {}
    for name, case in pc.CASES.items():
        r = pc.oracle_run(case, po.reference())
        assert r["begin"] == 0 and r["rhs_code"] == 0 and r["run"] == 0 and r["diag"] == 0, name
        for k in ["rate", "rhs", "H", "T", "phi"]:
            data[f"{name}_{k}"] = r[k]
        data[f"{name}_scalars"] = np.array([r["limit"], r["bflux"]])
        data[f"{name}_rows"] = np.array([[row[f] for f in ROW_FIELDS] for row in [r["first"]] + r["rows"]])
    np.savez_compressed(os.path.join(HERE, "preheat_golden.npz"), **data)
    print("preheat_golden.npz:", len(data), "arrays")


def quads_golden():
    """The reference-backed transport on perturbed-quadrilateral and
    sine-stretched meshes (src/core/mesh.cpp:27-55): one RHS with the limiter
    factors, and 10 SSPRK3 steps."""
    import quad_cases as qc
    data = {}
    for name in qc.QUAD_CASES:
        t, xy, _, _ = qc.quad_oracle(name, po.reference())
        code, r = t.rhs()
        assert code == 0, (name, code)
        code, thH, thC = t.limiter()
        assert code == 0
        for k in ["rhsH", "rhsC", "T", "phi", "rate"]:
            data[f"{name}_rhs_{k}"] = r[k]
        data[f"{name}_rhs_totals"] = np.array([r["boundaryH"], r["boundaryC"], r["maxRate"], r["divergence"]])
        data[f"{name}_thetaH"], data[f"{name}_thetaC"] = thH, thC
        data[f"{name}_xy"] = xy
        t, _, _, _ = qc.quad_oracle(name, po.reference())
        code, reps = t.step(10)
        assert code == 0, (name, code)
        data[f"{name}_rk3_10"] = np.stack(t.get_state())
        data[f"{name}_rk3_10_dt"] = np.array([x["dt"] for x in reps])
        data[f"{name}_rk3_10_retries"] = np.array([x["retries"] for x in reps])
    np.savez_compressed(os.path.join(HERE, "quads_golden.npz"), **data)
    print("quads_golden.npz:", len(data), "arrays")


if __name__ == "__main__":
    if not po.reference_available():
        sys.exit("reference build missing: run `make -C oracle ref` where the reference is mounted")
    which = sys.argv[1:] or ["phase", "transport", "preheat", "quads"]
    if "phase" in which:
        phase_golden()
    if "transport" in which:
        transport_golden()
    if "preheat" in which:
        preheat_golden()
    if "quads" in which:
        quads_golden()

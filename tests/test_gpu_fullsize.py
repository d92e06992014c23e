"""GPU parity at the full size of the headline workload: 1280x2560 uniform
quads, the bench's seeded construction (seed 1), SSPRK3 at CFL 0.4.

Compared cell by cell, |x - ref| / max(|ref|, 1e-3 max|ref|), at 1e-12:
the limiter factors theta_H, theta_C of the initial state; one stage L(U^n)
(T, phi, rate per cell; rhsH, rhsC against their infinity norm; the stage
totals); one accepted SSPRK3 step (dt, retries, H, C, T, phi).

Two stencil-table conventions exist for a uniform mesh. The reference builds
every cell's tables from that cell's own rounded vertex coordinates
(TensorStencilPoly::Initialize per cell, src/mlweno/tensorstencilpoly.cpp:
146-231). The headline path builds one table set per mesh (every cell of a
uniform mesh has the same stencil geometry up to that rounding); the
general-quad path (the same mesh given as vertices) builds per-cell tables
on the GPU as the reference does. Three comparisons run: headline path vs
the restated oracle with one table set per mesh (the same convention),
vertex path vs the per-cell-table oracle (the reference build), headline
path vs the per-cell-table oracle.

Every stage quantity and the step (rhsH, rhsC, rate, T, the stage totals,
dt, retries, H, C, T after the step) is held to 1e-12 in all three.

The limiter factors theta_H, theta_C and the fractions phi (stage and after
the step) are ratios whose per-cell relative error is the rounding of their
inputs times a condition number that is large in a few of the 3.3M cells:
theta = (bound - mean) / (extreme - mean) where the reconstruction barely
overshoots, phi just above the solidus. The reference's algorithm shows it
itself: the two oracles, which differ only by the rounding of stencil-table
entries (a few ulp), are up to 7e-12 (theta_H), 1e-11 (theta_C) and 5e-12
(phi) apart per cell at this size, and the same restatement evaluated with
double instead of long double intermediates moves theta by up to 8e-13. The
GPU's FP64 evaluation is another such rounding. These four are held to
1e-12 plus twice the distance between the two oracles measured in the same
run (the per-cell-table convention's own spread), and, cell by cell, the
cells above 1e-12 must be few (at most 0.1 %) and, 95 % of them or more,
cells where the two conventions of the reference differ by more than 1e-14.

The reference build needs about 23 KB of host memory per cell; where the
host has less free memory, the per-cell-table oracle is the restated one
(bit for bit the reference build on every golden case).
"""
import os

import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * max(np.max(np.abs(b)), 1e-300))))


def per_cell(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * max(np.max(np.abs(b)), 1e-300))


def rel_inf(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def host_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def gpu_run(w, vertices=None):
    from mantlepar_b200.transport import Transport, TransportConfig
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3), vertices=vertices)
    t.set_face_velocity(*(sy.face_velocity(w) if vertices is None else sy.face_velocity_quads(w, vertices)))
    t.set_state(*sy.initial_state(w))
    th = t.limiter()
    r = t.rhs()
    _, reps = t.step(1)
    st = t.get_state()
    t.close()
    return dict(th=th, rhs=r, rep=reps[0], st=st)


def oracle_run(w, lib, uniform):
    from oracle import pyoracle as po
    o = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=3, threads=os.cpu_count() or 1,
                           uniform_tables=uniform)
    o.set_face_velocity(*sy.face_velocity(w))
    o.set_state(*sy.initial_state(w))
    code, a, b = o.limiter()
    assert code == 0
    code, r = o.rhs()
    assert code == 0
    code, reps = o.step(1)
    assert code == 0
    st = o.get_state()
    o.close()
    return dict(th=(a, b), rhs=r, rep=reps[0], st=st)


def errors(g, o):
    e = {"thetaH": rel(g["th"][0], o["th"][0]), "thetaC": rel(g["th"][1], o["th"][1])}
    for k in ("T", "phi", "rate"):
        e[k] = rel(g["rhs"][k], o["rhs"][k])
    for k in ("rhsH", "rhsC"):
        e[k] = rel_inf(g["rhs"][k], o["rhs"][k])
    e["maxRate"] = abs(g["rhs"]["maxRate"] - o["rhs"]["maxRate"]) / o["rhs"]["maxRate"]
    e["boundaryH"] = abs(g["rhs"]["boundaryH"] - o["rhs"]["boundaryH"]) / max(1.0, abs(o["rhs"]["boundaryH"]))
    e["dt"] = abs(g["rep"]["dt"] - o["rep"]["dt"]) / o["rep"]["dt"]
    assert g["rep"]["retries"] == o["rep"]["retries"]
    for name, a, b in zip(("H", "C", "T1", "phi1"), g["st"], o["st"]):
        e[name] = rel(a, b)
    return e


def show(label, e):
    print(label, {k: f"{v:.2e}" for k, v in e.items()})


def test_headline_workload_against_the_oracles(cuda_lib):
    from oracle import pyoracle as po
    w = sy.Workload(nx=1280, ny=2560)
    g = gpu_run(w)
    gq = gpu_run(w, vertices=sy.quad_vertices(w, sy.MESH_RECTANGULAR))
    # Same table convention: the restated oracle with one table set per mesh.
    o_uni = oracle_run(w, po.restated(), True)
    e_uni = errors(g, o_uni)
    show("headline path vs restated oracle (one table set per mesh):", e_uni)
    # Per-cell tables: the reference build where the host has room for it.
    use_ref = po.reference_available() and host_available() > 1.5 * 23e3 * w.cells
    o_cell = oracle_run(w, po.reference() if use_ref else po.restated(), False)
    label = "reference build" if use_ref else "restated oracle (per-cell tables)"
    e_vtx = errors(gq, o_cell)
    show(f"vertex path vs {label}:", e_vtx)
    gap = errors(o_uni, o_cell)
    show(f"restated oracle (one table set) vs {label}:", gap)
    e_cell = errors(g, o_cell)
    show(f"headline path vs {label}:", e_cell)
    fractions = ("thetaH", "thetaC", "phi", "phi1")
    for e in (e_uni, e_vtx, e_cell):
        for k, v in e.items():
            bound = RTOL if k not in fractions else 2 * gap[k] + RTOL
            assert v <= bound, (k, v, bound)
    # Cell by cell: the few cells where the headline path moves a ratio by
    # more than 1e-12 (measured: 0.02-0.08 % of the cells) are, all but a
    # handful, cells where the reference's own value moves with the rounding
    # of its stencil tables (the two conventions differ there by > 1e-14).
    pick = {"thetaH": lambda r: r["th"][0], "thetaC": lambda r: r["th"][1],
            "phi": lambda r: r["rhs"]["phi"], "phi1": lambda r: r["st"][3]}
    for k in fractions:
        gv, uv, cv = pick[k](g), pick[k](o_uni), pick[k](o_cell)
        e_g = per_cell(gv, uv)
        big = e_g > RTOL
        sensitive = per_cell(uv, cv)[big] > 1e-14
        print(f"{k}: {int(big.sum())} cells above 1e-12, {int(sensitive.sum())} of them table-sensitive")
        assert big.mean() <= 1e-3, (k, big.mean())
        assert sensitive.mean() >= 0.95 if big.any() else True, (k, sensitive.mean())

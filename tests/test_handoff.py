"""Handoff files: cellH1.dat / cellC1.dat + transport_state.json written as the
reference writes them (initialization.cpp:645-680,823-840) and validated on
import as LoadPreheatState does (evolve.cpp:54-125); evolution_history.csv
columns of evolve.cpp:443."""
import json
import os

import numpy as np
import pytest

from mantlepar_b200 import handoff as ho
from mantlepar_b200 import synthetic as sy
from oracle import pyoracle as po

W = sy.Workload(nx=12, ny=9, seed=4)
DERIVED = {"h0": 1.2e6, "l0": 316227.7660168379, "t0": 6324555320.336759}


def state():
    return sy.initial_state(W)


def test_round_trip_is_exact(tmp_path):
    H, C = state()
    mesh = ho.MeshInfo.of(W)
    ho.write_state(str(tmp_path), mesh, H, C, 0.0123, 17, DERIVED)
    H2, C2, t = ho.read_state(str(tmp_path), mesh, DERIVED, Xe=0.5)
    assert np.array_equal(H2, H) and np.array_equal(C2, C) and t == 0.0123
    lines = open(tmp_path / "cellH1.dat").read().splitlines()
    assert len(lines) == W.ny and all(len(l.split(" ")) == W.nx for l in lines)
    assert float(lines[1].split(" ")[2]) == H[1 * W.nx + 2]          # natural order j*nx + i
    m = json.load(open(tmp_path / "transport_state.json"))
    assert m["schema_version"] == 1 and m["status"] == "complete" and m["accepted_steps"] == 17
    assert m["mesh"]["nx"] == W.nx and m["H"] == {"file": "cellH1.dat", "units": "h/(cp*dT)"}
    assert not any(f.endswith(".tmp") for f in os.listdir(tmp_path))


@pytest.mark.parametrize("edit,msg", [
    (lambda m: m.update(status="incomplete"), "complete schema 1"),
    (lambda m: m.update(ordering="i*ny+j"), "representation/order"),
    (lambda m: m["C"].update(units="percent"), "units"),
    (lambda m: m["mesh"].update(nx=13), "mesh does not match"),
    (lambda m: m["mesh"]["domain"].__setitem__(1, 0.6), "domain"),
    (lambda m: m["scales"].update(time_s=1.0), "scales"),
    (lambda m: m.update(time=float("nan")), "Nonfinite"),
])
def test_manifest_checks(tmp_path, edit, msg):
    H, C = state()
    mesh = ho.MeshInfo.of(W)
    ho.write_state(str(tmp_path), mesh, H, C, 0.0, 0, DERIVED)
    p = tmp_path / "transport_state.json"
    m = json.load(open(p))
    edit(m)
    p.write_text(json.dumps(m))
    with pytest.raises(ho.HandoffError, match=msg):
        ho.read_state(str(tmp_path), mesh, DERIVED, Xe=0.5)


@pytest.mark.parametrize("field,values,msg", [
    ("cellC1.dat", lambda C: np.where(np.arange(C.size) == 5, 0.6, C), "Inadmissible"),
    ("cellH1.dat", lambda H: np.where(np.arange(H.size) == 3, -1.0, H), "Inadmissible"),
    ("cellH1.dat", lambda H: np.append(H, 1.0), "Extra entries"),
    ("cellC1.dat", lambda C: C[:-1], "Incomplete"),
])
def test_matrix_checks(tmp_path, field, values, msg):
    H, C = state()
    mesh = ho.MeshInfo.of(W)
    ho.write_state(str(tmp_path), mesh, H, C, 0.0, 0, DERIVED)
    a = H if field == "cellH1.dat" else C
    (tmp_path / field).write_text(" ".join(format(v, ".17g") for v in values(a)) + "\n")
    with pytest.raises(ho.HandoffError, match=msg):
        ho.read_state(str(tmp_path), mesh, DERIVED, Xe=0.5)


def test_history_rows_from_oracle_steps(tmp_path):
    t = po.TransportOracle(sy.material_s(), W, integrator=3)
    vs, ud = sy.face_velocity(W)
    H, C = state()
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    mesh = ho.MeshInfo.of(W)
    path = str(tmp_path / "evolution_history.csv")
    with ho.HistoryWriter(path, mesh, DERIVED) as hw:
        _, _, _, phi = t.get_state()
        hw.row(0, 0.0, H, C, phi)
        for k in range(3):
            code, (r,) = t.step(1)
            assert code == 0
            h, c, _, phi = t.get_state()
            hw.row(k + 1, r["time"], h, c, phi, r, dt=r["dt"], courant=r["courant"], retries=r["retries"])
    rows = ho.read_history(path)
    assert open(path).readline().strip() == ho.HISTORY_COLUMNS
    assert [r["step"] for r in rows] == [0, 1, 2, 3]
    assert rows[0]["dt"] == 0.0 and rows[3]["courant"] <= 0.4 * (1 + 1e-12)
    assert abs(rows[3]["H_integral"] - r["H_integral"]) <= 1e-13 * abs(r["H_integral"])

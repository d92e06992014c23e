"""The C++ coupled-transport layer (include/mantle/couple/coupled_transport.h):
AdvancePhaseCoupled and RHS through tests/cpp/run_coupled.cpp agree bit for
bit with the same solve through the C ABI from Python, and with the oracle to
1e-11; time.end, the fixed control and time.maximumSteps behave as the
reference's Run (src/couple/evolve.cpp:449-483)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from mantlepar_b200 import synthetic as sy

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(cuda_lib, tmp_path_factory):
    from mantlepar_b200 import build
    build.build_host()
    exe = str(tmp_path_factory.mktemp("cpp") / "run_coupled")
    cxx = os.environ.get("CXX") or shutil.which("g++")
    pkg = os.path.join(ROOT, "mantlepar_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "run_coupled.cpp"), "-L", pkg,
                    "-l:libmantle_b200_host.so", "-l:libmantlepar_b200.so", f"-Wl,-rpath,{pkg}", "-o", exe],
                   check=True)
    return exe


def run(driver, tmp_path, w, t_end, control, dt0, integ, max_steps=100000):
    H, C = sy.initial_state(w)
    vs, ud = sy.face_velocity(w)
    head = np.array([w.nx, w.ny, w.x0, w.x1, w.y0, w.y1, t_end, control, dt0, w.cfl, integ, max_steps], float)
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    np.concatenate([head, H, C, np.ravel(vs), np.ravel(ud)]).tofile(inp)
    subprocess.run([driver, inp, out], check=True, capture_output=True, text=True, timeout=300)
    d = np.fromfile(out)
    n = w.cells
    st, rs, time, acc, ns = d[:5]
    o = 5
    rH, rC = d[o:o + n], d[o + n:o + 2 * n]
    o += 2 * n
    maxrate = d[o]
    o += 1
    state = d[o:o + 4 * n].reshape(4, n)
    o += 4 * n
    hist = d[o:o + 3 * int(ns)].reshape(-1, 3)
    return dict(status=int(st), rhs_status=int(rs), time=time, accepted=int(acc), rhsH=rH, rhsC=rC,
                maxRate=maxrate, state=state, hist=hist)


def rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * np.max(np.abs(b))))


@pytest.mark.parametrize("control,dt0", [(0, 1e30), (1, 2e-4)], ids=["cfl", "fixed"])
def test_advance_phase_coupled_matches_c_abi_and_oracle(driver, tmp_path, control, dt0):
    from oracle import pyoracle as po
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=20, ny=20)
    t_end = 0.0071
    got = run(driver, tmp_path, w, t_end, control, dt0, 3)
    assert got["status"] == 0 and got["rhs_status"] == 0
    assert got["time"] == t_end
    # the same solve through the C ABI from Python
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3, dt_initial=dt0))
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    r = t.rhs()
    assert np.array_equal(got["rhsH"], r["rhsH"]) and np.array_equal(got["rhsC"], r["rhsC"])
    assert got["maxRate"] == r["maxRate"]
    t.set_time_control(control, t_end)
    _, reps = t.step(200)
    taken = [x for x in reps if x["dt"] > 0]
    assert got["accepted"] == len(taken)
    assert np.array_equal(got["hist"][:, 0], [x["dt"] for x in taken])
    assert np.array_equal(got["hist"][:, 1], [x["retries"] for x in taken])
    assert np.array_equal(got["state"], np.stack(t.get_state()))
    # the oracle
    o = po.TransportOracle(sy.material_s(), w, integrator=3, dt_initial=dt0)
    o.set_face_velocity(vs, ud)
    o.set_state(H, C)
    o.set_time_control(control, t_end)
    code, _ = o.step(200)
    assert code == 0
    ref = np.stack(o.get_state())
    for k in range(4):
        assert rel(got["state"][k], ref[k]) <= 1e-11, k


def test_maximum_steps_stops_with_not_converged(driver, tmp_path):
    w = sy.Workload(nx=20, ny=20)
    got = run(driver, tmp_path, w, 1.0, 0, 1e30, 2, max_steps=3)
    assert got["status"] == 91 and got["accepted"] == 3 and len(got["hist"]) == 3


@pytest.fixture(scope="module")
def preheat_driver(cuda_lib, tmp_path_factory):
    from mantlepar_b200 import build
    build.build_host()
    exe = str(tmp_path_factory.mktemp("cpp") / "run_preheat")
    cxx = os.environ.get("CXX") or shutil.which("g++")
    pkg = os.path.join(ROOT, "mantlepar_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "run_preheat.cpp"), "-L", pkg,
                    "-l:libmantle_b200_host.so", "-l:libmantlepar_b200.so", f"-Wl,-rpath,{pkg}", "-o", exe],
                   check=True)
    return exe


@pytest.mark.parametrize("name", ["through_diffusion", "global_fixed", "quad_through"])
def test_advance_legacy_preheat_matches_reference(preheat_driver, tmp_path, name):
    """AdvanceLegacyPreheat and WritePreheatHistory (src/couple/preheat.cpp:
    235-312) through the C++ layer, on uniform and perturbed meshes: rows,
    final H, T and phi within 1e-12 of the reference-backed golden run; the
    CSV holds the reference's columns."""
    import preheat_cases as pc
    from mantlepar_b200.preheat import HISTORY_COLUMNS
    case = pc.CASES[name]
    w = case.w
    H, C = case.state()
    head = np.array([w.nx, w.ny, w.x0, w.x1, w.y0, w.y1, case.end, case.control, case.dt_initial, case.dt_min,
                     case.dt_max, case.cfl, case.max_steps, case.kappa, *case.thermal_type, *case.thermal_value,
                     case.H_policy, case.inflow_H, case.lf_global, case.lf_global_speed, case.pressure_model,
                     case.surface_y, 0.0 if case.family == 0 else 1.0, 0.0], float)
    assert head.size == 30
    inp, out, csv = str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), str(tmp_path / "preheat_history.csv")
    xy = case.vertices()
    np.concatenate([head, H, C, np.ravel(case.velocity())] + ([] if xy is None else [xy])).tofile(inp)
    subprocess.run([preheat_driver, inp, out, csv], check=True, capture_output=True, text=True, timeout=300)
    d = np.fromfile(out)
    n = w.cells
    st, time, acc, nrows = d[:4]
    assert int(st) == 0 and time == case.end
    Hf, T, phi = d[4:4 + n], d[4 + n:4 + 2 * n], d[4 + 2 * n:4 + 3 * n]
    rows = d[4 + 3 * n:4 + 3 * n + 9 * int(nrows)].reshape(-1, 9)
    rep = d[4 + 3 * n + 9 * int(nrows):]
    G = np.load(os.path.join(ROOT, "tests", "golden", "preheat_golden.npz"))
    ref = G[f"{name}_rows"]
    assert rows.shape == ref.shape and int(acc) == int(ref[-1][0])
    assert np.array_equal(rows[:, 0], ref[:, 0])
    assert np.max(np.abs(rows[:, 1:7] - ref[:, 1:7]) / np.maximum(np.abs(ref[:, 1:7]), 1e-300)) <= 1e-12
    assert rel(Hf, G[f"{name}_H"]) <= 1e-12 and rel(T, G[f"{name}_T"]) <= 1e-12
    assert rep[1] == case.end and abs(rep[4] - ref[-1][4]) <= 1e-12 * abs(ref[-1][4])
    lines = open(csv).read().splitlines()
    assert lines[0] == HISTORY_COLUMNS and len(lines) == 1 + ref.shape[0]
    last = [float(x) for x in lines[-1].split(",")]
    assert int(last[0]) == int(ref[-1][0]) and last[1] == rows[-1][1] and last[6] == rows[-1][4]
